// The context entry points of the C ABI: open/close, errors, cancel flag, progress.
#include "kg_internal.cuh"

namespace kg {
std::atomic<uint64_t> g_launches{0};
std::atomic<uint64_t> g_allocs_left{UINT64_MAX};

cudaMemPool_t device_pool(int device) {
  static std::mutex mu;
  static std::vector<cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  if ((size_t)device >= pools.size()) pools.resize((size_t)device + 1, nullptr);
  if (!pools[device]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    KG_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t threshold = UINT64_MAX;
    KG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    pools[device] = pool;
  }
  return pools[device];
}

thread_local bool g_stage_pageable = false;

namespace {

// Page-locked staging for pageable host sources: two 16 MB halves and an event each, per
// device (events belong to a device), kept on a free list for the process's lifetime.
constexpr size_t kStageBytes = 16u << 20;
struct Staging {
  void* half[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
};
std::mutex g_stage_mu;
std::vector<std::vector<Staging*>> g_stage_free;

Staging* take_staging(int device) {
  {
    std::lock_guard<std::mutex> lock(g_stage_mu);
    if ((size_t)device < g_stage_free.size() && !g_stage_free[device].empty()) {
      Staging* st = g_stage_free[device].back();
      g_stage_free[device].pop_back();
      return st;
    }
  }
  auto st = std::make_unique<Staging>();
  for (int b = 0; b < 2; ++b) {
    KG_CUDA(cudaHostAlloc(&st->half[b], kStageBytes, cudaHostAllocPortable));
    KG_CUDA(cudaEventCreateWithFlags(&st->done[b], cudaEventDisableTiming));
  }
  return st.release();
}

void give_staging(int device, Staging* st) {
  std::lock_guard<std::mutex> lock(g_stage_mu);
  if ((size_t)device >= g_stage_free.size()) g_stage_free.resize((size_t)device + 1);
  g_stage_free[device].push_back(st);
}

}  // namespace

void staged_copy_to_device(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
  int device = 0;
  KG_CUDA(cudaGetDevice(&device));
  Staging* st = take_staging(device);
  bool used[2] = {false, false};
  try {
    size_t i = 0;
    for (size_t off = 0; off < bytes; off += kStageBytes, ++i) {
      const int b = (int)(i & 1);
      const size_t n = std::min(kStageBytes, bytes - off);
      // The half's previous copy has read it before the host overwrites it.
      if (used[b]) KG_CUDA(cudaEventSynchronize(st->done[b]));
      std::memcpy(st->half[b], (const char*)src + off, n);
      KG_CUDA(cudaMemcpyAsync((char*)dst + off, st->half[b], n, cudaMemcpyHostToDevice, stream));
      KG_CUDA(cudaEventRecord(st->done[b], stream));
      used[b] = true;
    }
    for (int b = 0; b < 2; ++b)
      if (used[b]) KG_CUDA(cudaEventSynchronize(st->done[b]));
  } catch (...) {
    // Wait (unchecked) for copies already queued before the halves go back.
    for (int b = 0; b < 2; ++b)
      if (used[b]) cudaEventSynchronize(st->done[b]);
    give_staging(device, st);
    throw;
  }
  give_staging(device, st);
}

std::string& last_error() {
  thread_local std::string message;
  return message;
}

void trace_slow_alloc(size_t bytes, double ms) {
  int device = 0;
  uint64_t reserved = 0, used = 0;
  size_t free_b = 0, total_b = 0;
  if (cudaGetDevice(&device) == cudaSuccess) {
    cudaMemPool_t pool = device_pool(device);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
  }
  cudaMemGetInfo(&free_b, &total_b);
  std::fprintf(stderr,
               "[kyto_gpu trace] slow allocation: %.3f GB in %.1f ms (pool reserved %.2f GB, "
               "used %.2f GB; device free %.2f GB)\n",
               bytes / 1e9, ms, reserved / 1e9, used / 1e9, free_b / 1e9);
}
}  // namespace kg

extern "C" {

kg_status kg_open(int device, kg_ctx** out) {
  return kg::guarded([&] {
    if (!out) kg::fail(KG_ERR_INVALID, "kg_open: out is NULL");
    *out = nullptr;
    int n = 0;
    KG_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n)
      kg::fail(KG_ERR_INVALID, "kg_open: device " + std::to_string(device) +
                                   " does not exist (" + std::to_string(n) + " found)");
    KG_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop{};
    KG_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
      kg::fail(KG_ERR_INVALID, std::string("kg_open: ") + prop.name +
                                   " is not a Blackwell (sm_100a) device");
    auto* ctx = new kg_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    try {
      KG_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
      KG_CUBLAS(cublasCreate(&ctx->cublas));
      KG_CUSOLVER(cusolverDnCreate(&ctx->cusolver));
      // The library's own pool on this device (memory it frees stays there between
      // calls; the device's default pool is left as the process set it).
      kg::device_pool(device);
    } catch (...) {
      if (ctx->cusolver) cusolverDnDestroy(ctx->cusolver);
      if (ctx->cublas) cublasDestroy(ctx->cublas);
      if (ctx->stream) cudaStreamDestroy(ctx->stream);
      delete ctx;
      throw;
    }
    *out = ctx;
  });
}

void kg_close(kg_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->knn_ws.reset();
  cudaStreamSynchronize(ctx->stream);
  for (const kg_ctx::SessionRes& r : ctx->free_res) {
    cudaStreamSynchronize(r.stream);
    cusolverDnDestroy(r.cusolver);
    cublasDestroy(r.cublas);
    cudaStreamDestroy(r.stream);
  }
  if (ctx->cusolver) cusolverDnDestroy(ctx->cusolver);
  if (ctx->cublas) cublasDestroy(ctx->cublas);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

size_t kg_last_error(const kg_ctx*, char* buf, size_t len) {
  const std::string& m = kg::last_error();
  if (buf && len) {
    size_t n = m.size() < len - 1 ? m.size() : len - 1;
    std::memcpy(buf, m.data(), n);
    buf[n] = '\0';
  }
  return m.size();
}

kg_status kg_set_cancel_flag(kg_ctx* ctx, const volatile int32_t* flag) {
  return kg::guarded([&] {
    if (!ctx) kg::fail(KG_ERR_INVALID, "kg_set_cancel_flag: ctx is NULL");
    ctx->cancel = flag;
  });
}

kg_status kg_set_wait_limit(kg_ctx* ctx, double seconds) {
  return kg::guarded([&] {
    if (!ctx) kg::fail(KG_ERR_INVALID, "kg_set_wait_limit: ctx is NULL");
    if (!(seconds > 0.0)) kg::fail(KG_ERR_INVALID, "kg_set_wait_limit: seconds must be > 0");
    ctx->wait_limit_s = seconds;
  });
}

kg_status kg_reserve(kg_ctx* ctx, uint64_t bytes) {
  return kg::guarded([&] {
    if (!ctx) kg::fail(KG_ERR_INVALID, "kg_reserve: ctx is NULL");
    if (!bytes) return;
    KG_CUDA(cudaSetDevice(ctx->device));
    // The library pool's release threshold is the maximum: a freed block stays reserved.
    void* p = nullptr;
    KG_CUDA(cudaMallocFromPoolAsync(&p, bytes, kg::device_pool(ctx->device), ctx->stream));
    KG_CUDA(cudaFreeAsync(p, ctx->stream));
    KG_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

kg_status kg_progress(const kg_ctx* ctx, uint64_t* done, uint64_t* total) {
  return kg::guarded([&] {
    if (!ctx) kg::fail(KG_ERR_INVALID, "kg_progress: ctx is NULL");
    if (done) *done = ctx->done.load();
    if (total) *total = ctx->total.load();
  });
}

kg_status kg_diag_pool_usage(int device, uint64_t* reserved, uint64_t* used,
                             uint64_t* used_high, int32_t reset_high) {
  return kg::guarded([&] {
    int n = 0;
    KG_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) kg::fail(KG_ERR_INVALID, "kg_diag_pool_usage: no such device");
    cudaMemPool_t pool = kg::device_pool(device);
    uint64_t v = 0;
    if (reserved) KG_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, reserved));
    if (used) KG_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, used));
    if (used_high) KG_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, used_high));
    if (reset_high) KG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &v));
  });
}

kg_status kg_diag_fail_allocations(uint64_t after) {
  return kg::guarded([&] { kg::g_allocs_left.store(after); });
}

kg_status kg_diag_kernel_launches(uint64_t* count) {
  return kg::guarded([&] {
    if (!count) kg::fail(KG_ERR_INVALID, "kg_diag_kernel_launches: count is NULL");
    *count = kg::g_launches.load();
  });
}

}  // extern "C"
