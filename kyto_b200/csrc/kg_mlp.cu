// The learned partitioner's network (kg_mlp.cuh): forward, backward and Adam on the
// device. Every reduction runs in a fixed order (no float atomics), so training is
// bit-reproducible run to run.
#include "kg_mlp.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>

#include "kg_sm100.cuh"
#include "kg_tma.cuh"

namespace kg {

using namespace sm100;

namespace {

constexpr int kBM = 64, kBN = 64, kBK = 16;  // GEMM block tile
constexpr int kGemmThreads = 256;            // 16 x 16 threads, 4 x 4 outputs each

enum : int { kEpiStore = 0, kEpiBiasReluBf16 = 1, kEpiMaskRelu = 2, kEpiBias = 3 };

__device__ __forceinline__ float as_f32(float v) { return v; }
__device__ __forceinline__ float as_f32(__nv_bfloat16 v) { return __bfloat162float(v); }

// C (M x N, row stride ldc) = op(A) (M x K) . op(B) (K x N), f32 sums of bf16 or f32
// operands in k order per output (each output is one thread's running sum over the k
// tiles: a fixed order). A(m,k) = TA ? A[k*lda+m] : A[m*lda+k]; B(k,n) = TB ? B[n*ldb+k]
// : B[k*ldb+n]. Epilogues: store; + bias then ReLU rounded to bf16 into h (C keeps the
// pre-activation); C * (z > 0) (the ReLU's backward); + bias.
// Split over K (gridDim.z > 1, the store epilogue only): slice z sums k in
// [z * kslice, (z + 1) * kslice) and writes its M x N partial at C + z * M * N (row
// stride N); split_sum_kernel then adds the slices in order.
template <class TA, class TB, bool TRA, bool TRB, int EPI>
__global__ void __launch_bounds__(kGemmThreads)
gemm_kernel(int M, int N, int K, const TA* __restrict__ A, int lda, const TB* __restrict__ B,
            int ldb, float* __restrict__ C, int ldc, const float* __restrict__ bias,
            __nv_bfloat16* __restrict__ h, int ldh, const float* __restrict__ z, int ldz,
            int kslice) {
  __shared__ float as[kBK][kBM + 4];
  __shared__ float bs[kBK][kBN + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int k_begin = (int)blockIdx.z * kslice, k_end = min(K, k_begin + kslice);
  if (gridDim.z > 1) {
    C += (size_t)blockIdx.z * M * N;
    ldc = N;
  }
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  for (int k0 = k_begin; k0 < k_end; k0 += kBK) {
    // 64 x 16 of A and 16 x 64 of B, 4 elements a thread each.
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = threadIdx.x + e * kGemmThreads;  // 0..1023
      int mm, kk;
      if (TRA) {  // consecutive threads along m
        mm = idx & 63;
        kk = idx >> 6;
      } else {    // consecutive threads along k
        kk = idx & 15;
        mm = idx >> 4;
      }
      const int gm = m0 + mm, gk = k0 + kk;
      float v = 0.0f;
      if (gm < M && gk < k_end) v = as_f32(TRA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk]);
      as[kk][mm] = v;
      int nn, kb;
      if (TRB) {
        kb = idx & 15;
        nn = idx >> 4;
      } else {
        nn = idx & 63;
        kb = idx >> 6;
      }
      const int gn = n0 + nn, gkb = k0 + kb;
      float w = 0.0f;
      if (gn < N && gkb < k_end) w = as_f32(TRB ? B[(size_t)gn * ldb + gkb] : B[(size_t)gkb * ldb + gn]);
      bs[kb][nn] = w;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = as[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + ty * 4 + i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx * 4 + j;
      if (gn >= N) continue;
      float v = acc[i][j];
      if (EPI == kEpiBiasReluBf16 || EPI == kEpiBias) v += bias[gn];
      if (EPI == kEpiMaskRelu) v = z[(size_t)gm * ldz + gn] > 0.0f ? v : 0.0f;
      C[(size_t)gm * ldc + gn] = v;
      if (EPI == kEpiBiasReluBf16) h[(size_t)gm * ldh + gn] = __float2bfloat16_rn(fmaxf(v, 0.0f));
    }
  }
}

// C (row stride ldc) = the sum of `splits` M x N slices (row stride N) in slice order.
__global__ void split_sum_kernel(const float* part, int splits, int M, int N, float* C, int ldc) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)M * N) return;
  float t = 0.0f;
  for (int z = 0; z < splits; ++z) t += part[(uint64_t)z * M * N + i];
  C[(i / N) * (uint64_t)ldc + i % N] = t;
}

template <class TA, class TB, bool TRA, bool TRB, int EPI>
void gemm(int M, int N, int K, const TA* A, int lda, const TB* B, int ldb, float* C, int ldc,
          cudaStream_t s, const float* bias = nullptr, __nv_bfloat16* h = nullptr, int ldh = 0,
          const float* z = nullptr, int ldz = 0) {
  if (M == 0 || N == 0) return;
  dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
  // A long K over few output tiles (the weight gradients: K = the batch's rows) is split
  // so that about two waves of CTAs run; the slices' partial sums are added in a fixed
  // order, so the result is the same run to run.
  int splits = 1;
  if (EPI == kEpiStore) {
    const int tiles = (int)(grid.x * grid.y);
    while (tiles * splits < 256 && K / (splits * 2) >= 4 * kBK) splits *= 2;
  }
  const int kslice = ((K + splits - 1) / splits + kBK - 1) / kBK * kBK;
  grid.z = splits;
  if (splits == 1) {
    gemm_kernel<TA, TB, TRA, TRB, EPI><<<grid, kGemmThreads, 0, s>>>(
        M, N, K, A, lda, B, ldb, C, ldc, bias, h, ldh, z, ldz, K);
    KG_LAUNCH_CHECK();
    return;
  }
  DeviceBuffer<float> part((size_t)splits * M * N, s);
  gemm_kernel<TA, TB, TRA, TRB, EPI><<<grid, kGemmThreads, 0, s>>>(
      M, N, K, A, lda, B, ldb, part.ptr, N, bias, h, ldh, z, ldz, kslice);
  KG_LAUNCH_CHECK();
  split_sum_kernel<<<blocks_for((uint64_t)M * N, 256), 256, 0, s>>>(part.ptr, splits, M, N, C, ldc);
  KG_LAUNCH_CHECK();
}

// x (rows x din, stride ldx) rounded to bf16, rows of ld0 >= din (zeros past din).
__global__ void to_bf16_rows_kernel(const float* x, uint64_t rows, uint32_t din, uint64_t ldx,
                                    uint32_t ld0, __nv_bfloat16* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= rows * ld0) return;
  uint64_t r = i / ld0, c = i % ld0;
  out[i] = __float2bfloat16_rn(c < din ? x[r * ldx + c] : 0.0f);
}

// ---------------------------------------------------------------- tensor-core layers --
//
// One layer's z = A W^T + b on the 5th-generation tensor cores: A (rows x K bf16, K a
// multiple of 64 up to 256) and W (N x K bf16, row-major: K-major like A), f32 sums in
// tensor memory. One CTA per 128-row x tn-column tile (tn = min(N, 256)), 128 threads:
// thread 0 loads every K block of both tiles by TMA (128-byte swizzle) and issues the
// MMAs (M = 128, N = tn, K = 16); then each thread reads its row from TMEM and writes
// z (f32) and, for a hidden layer, h = bf16(relu(z)).
constexpr int kTcRows = 128, kTcNMax = 256, kTcKMax = 256, kTcKBox = 64;

struct MlpTcSmem {
  uint8_t a[kTcKMax / kTcKBox][kTcRows * 128];  // K blocks of the rows' tile
  uint8_t b[kTcKMax / kTcKBox][kTcNMax * 128];  // K blocks of the weights' tile
  uint64_t full, done;
  uint32_t tmem_base;
  int abort;
};
constexpr size_t kMlpTcSmemBytes = sizeof(MlpTcSmem) + 1024;
static_assert(kMlpTcSmemBytes <= 227 * 1024, "MLP layer shared memory");

template <int EPI>
__global__ void __launch_bounds__(128, 1)
mlp_tc_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
              int M, int K, int tn, uint32_t idesc, const float* __restrict__ bias, float* z,
              int ldz, __nv_bfloat16* h, int ldh, int* error) {
  extern __shared__ uint8_t smem_raw[];
  MlpTcSmem& sm = *reinterpret_cast<MlpTcSmem*>(smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * kTcRows, n0 = blockIdx.x * tn;
  const int kb = K / kTcKBox;
  volatile int* abort = &sm.abort;
  if (threadIdx.x == 0) {
    mbar_init(&sm.full, 1);
    mbar_init(&sm.done, 1);
    sm.abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(&sm.tmem_base, kTcNMax);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;
  if (threadIdx.x == 0) {
    prefetch_tmap(&ta);
    prefetch_tmap(&tb);
    mbar_arrive_expect_tx(&sm.full, (uint32_t)kb * (uint32_t)(kTcRows + tn) * 128u);
    for (int j = 0; j < kb; ++j) {
      tma_load_2d(sm.a[j], &ta, &sm.full, j * kTcKBox, m0);
      tma_load_2d(sm.b[j], &tb, &sm.full, j * kTcKBox, n0);
    }
    if (mbar_wait(&sm.full, 0, abort)) {
      tc_fence_after();
      for (int j = 0; j < kb; ++j) {
        const uint32_t aa = smem_addr(sm.a[j]), bb = smem_addr(sm.b[j]);
#pragma unroll
        for (int kk = 0; kk < kTcKBox / 16; ++kk)
          mma_f16(tmem, desc_k_sw128(aa + kk * 32), desc_k_sw128(bb + kk * 32), idesc,
                  (j | kk) > 0);
      }
    } else {
      // The loads never all landed: let them finish (bounded) before the CTA leaves.
      for (uint32_t i = 0; i < kWaitPolls && !mbar_try_wait(&sm.full, 0); ++i) __nanosleep(64);
    }
    mma_commit(&sm.done);
  }
  __syncwarp();
  const bool ok = mbar_wait(&sm.done, 0, abort);
  tc_fence_after();
  __syncwarp();
  if (ok && !*abort) {
    const int row = m0 + warp * 32 + lane;
    for (int c = 0; c < tn / 32; ++c) {
      uint32_t r[32];
      tmem_ld_32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c * 32u, r);
      tmem_wait_ld();
      if (row >= M) continue;
      const int n = n0 + c * 32;
      float v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]) + bias[n + j];
      float4* zp = reinterpret_cast<float4*>(z + (size_t)row * ldz + n);
#pragma unroll
      for (int j = 0; j < 8; ++j)
        zp[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
      if (EPI == kEpiBiasReluBf16) {
        uint32_t packed[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const __nv_bfloat162 pr =
              __floats2bfloat162_rn(fmaxf(v[2 * j], 0.0f), fmaxf(v[2 * j + 1], 0.0f));
          packed[j] = *reinterpret_cast<const uint32_t*>(&pr);
        }
        uint4* hp = reinterpret_cast<uint4*>(h + (size_t)row * ldh + n);
#pragma unroll
        for (int j = 0; j < 4; ++j)
          hp[j] = make_uint4(packed[4 * j], packed[4 * j + 1], packed[4 * j + 2], packed[4 * j + 3]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (*abort && threadIdx.x == 0) atomicExch(error, 1);
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTcNMax);
  }
}

template <int EPI>
void mlp_tc_gemm(int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* W,
                 int ldw, const float* bias, float* z, int ldz, __nv_bfloat16* h, int ldh,
                 int* error, cudaStream_t s) {
  if (M == 0) return;
  const int tn = N < kTcNMax ? N : kTcNMax;
  if (K % kTcKBox || K > kTcKMax || tn % 32 || N % tn)
    fail(KG_ERR_INVALID, "MLP layer: shape outside the tensor-core tiles");
  static std::once_flag attr;
  std::call_once(attr, [] {
    KG_CUDA(cudaFuncSetAttribute(mlp_tc_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kMlpTcSmemBytes));
  });
  const CUtensorMap ta = tma_map_2d_16bit(A, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (uint64_t)K,
                                          (uint64_t)M, (uint64_t)lda * 2, kTcKBox, kTcRows);
  const CUtensorMap tb = tma_map_2d_16bit(W, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (uint64_t)K,
                                          (uint64_t)N, (uint64_t)ldw * 2, kTcKBox, (uint32_t)tn);
  const uint32_t idesc = idesc_f32acc(1u, kTcRows, (uint32_t)tn);
  dim3 grid((unsigned)(N / tn), (unsigned)((M + kTcRows - 1) / kTcRows));
  mlp_tc_kernel<EPI><<<grid, 128, kMlpTcSmemBytes, s>>>(ta, tb, M, K, tn, idesc, bias, z, ldz, h,
                                                        ldh, error);
  KG_LAUNCH_CHECK();
}

// W1 (hidden x din) as bf16 rows of 64 (zeros past din): the first layer's tensor-core
// operand.
__global__ void pad_w1_kernel(const float* w1, uint32_t hidden, uint32_t din, __nv_bfloat16* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)hidden * 64) return;
  const uint64_t r = i / 64, c = i % 64;
  out[i] = __float2bfloat16_rn(c < din ? w1[r * din + c] : 0.0f);
}

// One warp per row: p = softmax(z); dz = (p - t) / rows with t the share of each part
// among the row's L labels; row_loss = -(1/L) sum over labels of log p[label].
__global__ void softmax_xent_kernel(const float* z, uint32_t rows, uint32_t parts,
                                    const uint32_t* labels, uint32_t L, float* dz,
                                    float* row_loss) {
  const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (row >= rows) return;
  const float* zr = z + (uint64_t)row * parts;
  float m = -INFINITY;
  for (uint32_t p = lane; p < parts; p += 32) m = fmaxf(m, zr[p]);
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  float sum = 0.0f;
  for (uint32_t p = lane; p < parts; p += 32) sum += __expf(zr[p] - m);
  for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
  const float inv_rows = 1.0f / (float)rows, inv_sum = 1.0f / sum;
  float* dr = dz + (uint64_t)row * parts;
  for (uint32_t p = lane; p < parts; p += 32) dr[p] = __expf(zr[p] - m) * inv_sum * inv_rows;
  __syncwarp();
  if (lane == 0) {
    const float share = inv_rows / (float)L;
    const float log_sum = logf(sum);
    float loss = 0.0f;
    for (uint32_t j = 0; j < L; ++j) {
      const uint32_t p = labels[(uint64_t)row * L + j];
      dr[p] -= share;
      loss -= zr[p] - m - log_sum;
    }
    row_loss[row] = loss / (float)L;
  }
}

// out[c] = sum over rows of a[r * ld + c], 16 row classes per column summed in order,
// then the classes in order.
__global__ void __launch_bounds__(1024)
column_sums_kernel(const float* a, uint32_t rows, uint32_t cols, uint32_t ld, float* out) {
  __shared__ float part[16][64];
  const uint32_t c = blockIdx.x * 64 + (threadIdx.x & 63u), cls = threadIdx.x >> 6;
  float t = 0.0f;
  if (c < cols)
    for (uint32_t r = cls; r < rows; r += 16) t += a[(uint64_t)r * ld + c];
  part[cls][threadIdx.x & 63u] = t;
  __syncthreads();
  if (cls == 0 && c < cols) {
    float u = 0.0f;
    for (int k = 0; k < 16; ++k) u += part[k][threadIdx.x & 63u];
    out[c] = u;
  }
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, uint64_t n, float lr,
                            float b1, float b2, float c1, float c2, float eps) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void refresh_kernel(const float* p, uint64_t n, __nv_bfloat16* wb) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) wb[i] = __float2bfloat16_rn(p[i]);
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// He-uniform weights U(-sqrt(6/fan_in), sqrt(6/fan_in)) from a counter-based stream
// (SplitMix64 of seed and position); biases stay zero.
__global__ void init_kernel(float* p, uint64_t begin, uint64_t n, uint32_t fan_in,
                            uint64_t seed) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t bits = mix64(seed * 0x9E3779B97F4A7C15ull + begin + i + 1);
  const double u = (double)(bits >> 11) * 0x1p-53;  // [0, 1)
  const double lim = sqrt(6.0 / (double)fan_in);
  p[begin + i] = (float)((2.0 * u - 1.0) * lim);
}

// The top `probe` parts of each row's logits (ties to the lower part): one warp per
// row, `probe` rounds of a warp argmax. The confidence is their summed softmax at each
// temperature temps[t] (the logits times temps[t]): conf[t * conf_stride + row].
constexpr uint32_t kMaxTemps = 16;
__global__ void top_parts_kernel(const float* z, uint64_t rows, uint32_t parts, uint32_t probe,
                                 const float* temps, uint32_t n_temps, uint32_t* top,
                                 float* conf, uint64_t conf_stride, uint32_t n_mass,
                                 uint16_t* mass_part, float* mass_prob) {
  const uint64_t row = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (row >= rows) return;
  const float* zr = z + row * parts;
  float m = -INFINITY;
  for (uint32_t p = lane; p < parts; p += 32) m = fmaxf(m, zr[p]);
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  float sum0 = 0.0f;  // the first temperature's normaliser, for the kept probabilities
  if (n_mass) {
    for (uint32_t p = lane; p < parts; p += 32) sum0 += __expf(temps[0] * (zr[p] - m));
    for (int o = 16; o; o >>= 1) sum0 += __shfl_xor_sync(0xFFFFFFFFu, sum0, o);
  }
  float picked[kMaxTemps];
  for (uint32_t t = 0; t < n_temps; ++t) picked[t] = 0.0f;
  uint32_t prev_p = 0xFFFFFFFFu;
  float prev_v = INFINITY;
  const uint32_t rounds = max(probe, n_mass);
  for (uint32_t t = 0; t < rounds; ++t) {
    // The best (value, part) strictly after (prev_v, prev_p) in the order.
    float bv = -INFINITY;
    uint32_t bp = 0xFFFFFFFFu;
    for (uint32_t p = lane; p < parts; p += 32) {
      const float v = zr[p];
      const bool after = v < prev_v || (v == prev_v && p > prev_p);
      if (after && (v > bv || (v == bv && p < bp))) {
        bv = v;
        bp = p;
      }
    }
    for (int o = 16; o; o >>= 1) {
      const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
      const uint32_t op = __shfl_xor_sync(0xFFFFFFFFu, bp, o);
      if (ov > bv || (ov == bv && op < bp)) {
        bv = ov;
        bp = op;
      }
    }
    if (t < n_mass && lane == 0) {
      mass_part[row * n_mass + t] = (uint16_t)bp;
      mass_prob[row * n_mass + t] = __expf(temps[0] * (bv - m)) / sum0;
    }
    if (t < probe) {
      if (lane == 0) top[row * probe + t] = bp;
      for (uint32_t i = 0; i < n_temps; ++i) picked[i] += __expf(temps[i] * (bv - m));
    }
    prev_v = bv;
    prev_p = bp;
  }
  for (uint32_t i = 0; i < n_temps; ++i) {
    float sum = 0.0f;
    for (uint32_t p = lane; p < parts; p += 32) sum += __expf(temps[i] * (zr[p] - m));
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
    if (lane == 0) conf[i * conf_stride + row] = picked[i] / sum;
  }
}

}  // namespace

void MlpShape::layout() {
  uint64_t o = 0;
  auto take = [&](uint64_t n) {  // 8 elements: 16-byte aligned as bf16 too
    uint64_t at = o;
    o += (n + 7) & ~7ull;
    return at;
  };
  for (int l = 0; l < 3; ++l) {
    w_off[l] = take((uint64_t)out(l) * in(l));
    b_off[l] = take(out(l));
  }
  total = o;
}

void MlpBatch::alloc(const MlpShape& sh, uint32_t n, cudaStream_t s) {
  rows = n;
  h0.alloc((uint64_t)n * sh.h0_ld(), s);
  h1.alloc((uint64_t)n * sh.hidden, s);
  h2.alloc((uint64_t)n * sh.hidden, s);
  z1.alloc((uint64_t)n * sh.hidden, s);
  z2.alloc((uint64_t)n * sh.hidden, s);
  z3.alloc((uint64_t)n * sh.parts, s);
  dz3.alloc((uint64_t)n * sh.parts, s);
  dz2.alloc((uint64_t)n * sh.hidden, s);
  dz1.alloc((uint64_t)n * sh.hidden, s);
  row_loss.alloc(n, s);
}

void Mlp::init(uint32_t din, uint32_t hidden, uint32_t parts, uint64_t seed, cudaStream_t s) {
  sh.din = din;
  sh.hidden = hidden;
  sh.parts = parts;
  sh.layout();
  params.alloc(sh.total, s);
  params.zero();
  grads.alloc(sh.total, s);
  grads.zero();
  m1.alloc(sh.total, s);
  m1.zero();
  m2.alloc(sh.total, s);
  m2.zero();
  wb.alloc(sh.total, s);
  if (sh.tensor_cores()) w1p.alloc((uint64_t)sh.hidden * 64, s);
  tc_error.alloc(1, s);
  tc_error.zero();
  for (int l = 0; l < 3; ++l) {
    uint64_t nw = (uint64_t)sh.out(l) * sh.in(l);
    init_kernel<<<blocks_for(nw, 256), 256, 0, s>>>(params.ptr, sh.w_off[l], nw, sh.in(l), seed);
    KG_LAUNCH_CHECK();
  }
  step = 0;
  refresh(s);
}

__global__ void centre_init_kernel(float* p, MlpShape sh, const double* c, uint32_t K,
                                   uint32_t ldc, float beta) {
  const uint32_t din = sh.din, H = sh.hidden, P = sh.parts;
  const uint64_t n1 = 2ull * din * din, n2 = 2ull * din * H, n3 = (uint64_t)P * H;
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n1) {  // W1 rows 0..2din: +e_r, then -e_(r - din)
    const uint64_t r = i / din, j = i % din;
    p[sh.w_off[0] + r * din + j] = r < din ? (j == r ? 1.0f : 0.0f) : (j == r - din ? -1.0f : 0.0f);
    return;
  }
  i -= n1;
  if (i < n2) {  // W2 rows 0..2din: the identity on units 0..2din
    const uint64_t r = i / H, j = i % H;
    p[sh.w_off[1] + r * H + j] = j == r ? 1.0f : 0.0f;
    return;
  }
  i -= n2;
  if (i < n3) {  // W3: 2 beta c_j on relu(x), -2 beta c_j on relu(-x), 0 elsewhere
    const uint64_t r = i / H, j = i % H;
    float v = 0.0f;
    if (r < K && j < din) v = (float)(2.0 * beta * c[r * ldc + j]);
    else if (r < K && j < 2ull * din) v = (float)(-2.0 * beta * c[r * ldc + (j - din)]);
    p[sh.w_off[2] + r * H + j] = v;
    return;
  }
  i -= n3;
  if (i < P) {  // b3: -beta |c_j|^2 (a part without a centre: far below the others)
    double sq = 0.0;
    if (i < K)
      for (uint32_t j = 0; j < din; ++j) sq += c[i * ldc + j] * c[i * ldc + j];
    p[sh.b_off[2] + i] = i < K ? (float)(-beta * sq) : -1e4f;
  }
}

void Mlp::init_from_centres(const double* centres, uint32_t K, uint32_t ldc, float beta,
                            cudaStream_t s) {
  if (sh.hidden < 2 * sh.din) fail(KG_ERR_INVALID, "centre init: hidden below 2 x inputs");
  if (K > sh.parts) fail(KG_ERR_INVALID, "centre init: more centres than parts");
  const uint64_t total = 2ull * sh.din * sh.din + 2ull * sh.din * sh.hidden +
                         (uint64_t)sh.parts * sh.hidden + sh.parts;
  centre_init_kernel<<<blocks_for(total, 256), 256, 0, s>>>(params.ptr, sh, centres, K, ldc,
                                                            beta);
  KG_LAUNCH_CHECK();
  refresh(s);
}

void Mlp::set_params(const float* src, cudaStream_t s) {
  KG_CUDA(cudaMemcpyAsync(params.ptr, src, sh.total * 4, cudaMemcpyDefault, s));
  refresh(s);
}

void Mlp::refresh(cudaStream_t s) {
  refresh_kernel<<<blocks_for(sh.total, 256), 256, 0, s>>>(params.ptr, sh.total, wb.ptr);
  KG_LAUNCH_CHECK();
  if (sh.tensor_cores()) {
    pad_w1_kernel<<<blocks_for((uint64_t)sh.hidden * 64, 256), 256, 0, s>>>(
        params.ptr + sh.w_off[0], sh.hidden, sh.din, w1p.ptr);
    KG_LAUNCH_CHECK();
  }
}

void Mlp::check(cudaStream_t s) const {
  int h = 0;
  KG_CUDA(cudaMemcpyAsync(&h, tc_error.ptr, 4, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  if (h) fail(KG_ERR_TIMEOUT, "an MLP layer on the tensor cores gave up waiting on its loads");
}

void Mlp::forward(const float* x, uint64_t ldx, MlpBatch& b, cudaStream_t s) const {
  const int n = (int)b.rows, din = (int)sh.din, h = (int)sh.hidden, P = (int)sh.parts;
  const int ld0 = (int)sh.h0_ld();
  to_bf16_rows_kernel<<<blocks_for((uint64_t)n * ld0, 256), 256, 0, s>>>(x, n, din, ldx, ld0,
                                                                        b.h0.ptr);
  KG_LAUNCH_CHECK();
  const __nv_bfloat16* W = wb.ptr;
  const float* bias = params.ptr;
  if (sh.tensor_cores()) {
    mlp_tc_gemm<kEpiBiasReluBf16>(n, h, ld0, b.h0.ptr, ld0, w1p.ptr, ld0, bias + sh.b_off[0],
                                  b.z1.ptr, h, b.h1.ptr, h, tc_error.ptr, s);
    mlp_tc_gemm<kEpiBiasReluBf16>(n, h, h, b.h1.ptr, h, W + sh.w_off[1], h, bias + sh.b_off[1],
                                  b.z2.ptr, h, b.h2.ptr, h, tc_error.ptr, s);
    mlp_tc_gemm<kEpiBias>(n, P, h, b.h2.ptr, h, W + sh.w_off[2], h, bias + sh.b_off[2], b.z3.ptr,
                          P, nullptr, 0, tc_error.ptr, s);
    return;
  }
  // z = h W^T + b: W is out x in row-major, so B(k, n) = W[n * in + k].
  gemm<__nv_bfloat16, __nv_bfloat16, false, true, kEpiBiasReluBf16>(
      n, h, din, b.h0.ptr, ld0, W + sh.w_off[0], din, b.z1.ptr, h, s, bias + sh.b_off[0],
      b.h1.ptr, h);
  gemm<__nv_bfloat16, __nv_bfloat16, false, true, kEpiBiasReluBf16>(
      n, h, h, b.h1.ptr, h, W + sh.w_off[1], h, b.z2.ptr, h, s, bias + sh.b_off[1], b.h2.ptr, h);
  gemm<__nv_bfloat16, __nv_bfloat16, false, true, kEpiBias>(
      n, P, h, b.h2.ptr, h, W + sh.w_off[2], h, b.z3.ptr, P, s, bias + sh.b_off[2]);
}

void Mlp::backward(const uint32_t* labels, uint32_t L, MlpBatch& b, cudaStream_t s) {
  const int n = (int)b.rows, din = (int)sh.din, h = (int)sh.hidden, P = (int)sh.parts;
  softmax_xent_kernel<<<blocks_for((uint64_t)n * 32, 256), 256, 0, s>>>(
      b.z3.ptr, n, P, labels, L, b.dz3.ptr, b.row_loss.ptr);
  KG_LAUNCH_CHECK();
  const __nv_bfloat16* W = wb.ptr;
  float* G = grads.ptr;
  // Layer 3: dW3 = dz3^T h2 (P x h), db3 = column sums of dz3, dz2 = (dz3 W3) * (z2 > 0).
  gemm<float, __nv_bfloat16, true, false, kEpiStore>(P, h, n, b.dz3.ptr, P, b.h2.ptr, h,
                                                     G + sh.w_off[2], h, s);
  column_sums_kernel<<<(P + 63) / 64, 1024, 0, s>>>(b.dz3.ptr, n, P, P, G + sh.b_off[2]);
  KG_LAUNCH_CHECK();
  gemm<float, __nv_bfloat16, false, false, kEpiMaskRelu>(n, h, P, b.dz3.ptr, P, W + sh.w_off[2],
                                                         h, b.dz2.ptr, h, s, nullptr, nullptr, 0,
                                                         b.z2.ptr, h);
  // Layer 2.
  gemm<float, __nv_bfloat16, true, false, kEpiStore>(h, h, n, b.dz2.ptr, h, b.h1.ptr, h,
                                                     G + sh.w_off[1], h, s);
  column_sums_kernel<<<(h + 63) / 64, 1024, 0, s>>>(b.dz2.ptr, n, h, h, G + sh.b_off[1]);
  KG_LAUNCH_CHECK();
  gemm<float, __nv_bfloat16, false, false, kEpiMaskRelu>(n, h, h, b.dz2.ptr, h, W + sh.w_off[1],
                                                         h, b.dz1.ptr, h, s, nullptr, nullptr, 0,
                                                         b.z1.ptr, h);
  // Layer 1.
  gemm<float, __nv_bfloat16, true, false, kEpiStore>(h, din, n, b.dz1.ptr, h, b.h0.ptr,
                                                     (int)sh.h0_ld(), G + sh.w_off[0], din, s);
  column_sums_kernel<<<(h + 63) / 64, 1024, 0, s>>>(b.dz1.ptr, n, h, h, G + sh.b_off[0]);
  KG_LAUNCH_CHECK();
}

void Mlp::adam(float lr, cudaStream_t s) {
  ++step;
  const float c1 = 1.0f - (float)std::pow(0.9, (double)step);
  const float c2 = 1.0f - (float)std::pow(0.999, (double)step);
  adam_kernel<<<blocks_for(sh.total, 256), 256, 0, s>>>(params.ptr, grads.ptr, m1.ptr, m2.ptr,
                                                        sh.total, lr, 0.9f, 0.999f, c1, c2, 1e-8f);
  KG_LAUNCH_CHECK();
  refresh(s);
}

// The same selection for rows of at most 1,024 parts with the row held in registers
// (lane l: parts l, l + 32, ...): each lane keeps its best part not yet taken, a round
// takes the warp's best of those (ties to the lower part) and only the lane that gave it
// looks again. Parts, probabilities and sums come out in the same order and bits as
// top_parts_kernel's.
constexpr uint32_t kRegParts = 32;  // parts a lane holds
__device__ __forceinline__ uint32_t order_key(float v) {
  const uint32_t b = __float_as_uint(v);
  return b ^ ((b >> 31) ? 0xFFFFFFFFu : 0x80000000u);  // unsigned order = float order
}

__global__ void __launch_bounds__(256)
top_parts_reg_kernel(const float* z, uint64_t rows, uint32_t parts, uint32_t probe,
                     const float* temps, uint32_t n_temps, uint32_t* top, float* conf,
                     uint64_t conf_stride, uint32_t n_mass, uint16_t* mass_part,
                     float* mass_prob) {
  const uint64_t row = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (row >= rows) return;
  const float* zr = z + row * parts;
  float v[kRegParts];
#pragma unroll
  for (uint32_t j = 0; j < kRegParts; ++j) {
    const uint32_t p = lane + 32 * j;
    v[j] = p < parts ? zr[p] : -INFINITY;
  }
  float m = -INFINITY;
#pragma unroll
  for (uint32_t j = 0; j < kRegParts; ++j) m = fmaxf(m, v[j]);
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  auto lane_sum = [&](float t) {
    float sum = 0.0f;
#pragma unroll
    for (uint32_t j = 0; j < kRegParts; ++j)
      if (lane + 32 * j < parts) sum += __expf(t * (v[j] - m));
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
    return sum;
  };
  const float sum0 = n_mass ? lane_sum(temps[0]) : 0.0f;
  // The lane's four best parts not yet taken, best first (value, then the lower slot on
  // ties), kept sorted; refilled from every slot when they run out.
  uint32_t taken = 0;
  float cv[4];
  uint32_t cj[4];
  auto refill = [&]() {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      cv[i] = -INFINITY;
      cj[i] = 0xFFFFFFFFu;
    }
#pragma unroll
    for (uint32_t j = 0; j < kRegParts; ++j) {
      if (lane + 32 * j >= parts || ((taken >> j) & 1u)) continue;
      float x = v[j];
      uint32_t xj = j;
      // Insert (strictly greater moves ahead: an earlier slot stays ahead on ties).
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const bool ahead = cj[i] == 0xFFFFFFFFu || x > cv[i];
        const float tv = cv[i];
        const uint32_t tj = cj[i];
        cv[i] = ahead ? x : cv[i];
        cj[i] = ahead ? xj : cj[i];
        x = ahead ? tv : x;
        xj = ahead ? tj : xj;
      }
    }
  };
  refill();
  float picked[kMaxTemps];
#pragma unroll
  for (uint32_t t = 0; t < kMaxTemps; ++t) picked[t] = 0.0f;
  // Round t's part and value are kept by lane t % 32 (rounds 32..63 in the second pair).
  uint32_t my_part0 = 0u, my_part1 = 0u;
  float my_val0 = 0.0f, my_val1 = 0.0f;
  const uint32_t rounds = max(probe, n_mass);
  for (uint32_t t = 0; t < rounds; ++t) {
    // The warp's best: the largest value, then the lowest part among the lanes with it.
    const bool live = cj[0] != 0xFFFFFFFFu;
    const uint32_t key = live ? order_key(cv[0]) : 0u;
    const uint32_t kmax = __reduce_max_sync(0xFFFFFFFFu, key);
    const uint32_t mine = (live && key == kmax) ? lane + 32 * cj[0] : 0xFFFFFFFFu;
    const uint32_t bp = __reduce_min_sync(0xFFFFFFFFu, mine);
    const float bv = __shfl_sync(0xFFFFFFFFu, cv[0], bp & 31u);
    if ((t & 31u) == lane) {
      if (t < 32) {
        my_part0 = bp;
        my_val0 = bv;
      } else {
        my_part1 = bp;
        my_val1 = bv;
      }
    }
    if (t < probe) {
#pragma unroll
      for (uint32_t i = 0; i < kMaxTemps; ++i)
        if (i < n_temps) picked[i] += __expf(temps[i] * (bv - m));
    }
    if (bp % 32 == lane) {
      taken |= 1u << (bp / 32);
      cv[0] = cv[1];
      cj[0] = cj[1];
      cv[1] = cv[2];
      cj[1] = cj[2];
      cv[2] = cv[3];
      cj[2] = cj[3];
      cv[3] = -INFINITY;
      cj[3] = 0xFFFFFFFFu;
      if (cj[0] == 0xFFFFFFFFu) refill();
    }
  }
#pragma unroll
  for (uint32_t h = 0; h < 2; ++h) {
    const uint32_t t = lane + 32 * h;
    const uint32_t part = h ? my_part1 : my_part0;
    const float val = h ? my_val1 : my_val0;
    if (t < probe) top[row * probe + t] = part;
    if (t < n_mass) {
      mass_part[row * n_mass + t] = (uint16_t)part;
      mass_prob[row * n_mass + t] = __expf(temps[0] * (val - m)) / sum0;
    }
  }
#pragma unroll
  for (uint32_t i = 0; i < kMaxTemps; ++i) {
    if (i >= n_temps) break;
    const float sum = lane_sum(temps[i]);
    if (lane == 0) conf[i * conf_stride + row] = picked[i] / sum;
  }
}

void top_parts(const float* logits, uint64_t rows, uint32_t parts, uint32_t probe, uint32_t* top,
               float* confidence, uint64_t conf_stride, cudaStream_t s, const float* temps,
               uint32_t n_temps, uint32_t n_mass, uint16_t* mass_part, float* mass_prob) {
  if (n_temps < 1 || n_temps > kMaxTemps) fail(KG_ERR_INVALID, "top_parts: 1..16 temperatures");
  if (n_mass > parts || parts > 65536) fail(KG_ERR_INVALID, "top_parts: kept parts");
  if (parts <= 32 * kRegParts && std::max(probe, n_mass) <= parts) {
    top_parts_reg_kernel<<<blocks_for(rows * 32, 256), 256, 0, s>>>(
        logits, rows, parts, probe, temps, n_temps, top, confidence, conf_stride, n_mass,
        mass_part, mass_prob);
    KG_LAUNCH_CHECK();
    return;
  }
  top_parts_kernel<<<blocks_for(rows * 32, 256), 256, 0, s>>>(logits, rows, parts, probe, temps,
                                                             n_temps, top, confidence,
                                                             conf_stride, n_mass, mass_part,
                                                             mass_prob);
  KG_LAUNCH_CHECK();
}

}  // namespace kg
