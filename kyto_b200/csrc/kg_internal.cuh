// Internal helpers of libkyto_gpu.so: errors, the context, device buffers, bounded
// waits. Nothing here crosses the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <mutex>
#include <string>
#include <thread>
#include <utility>

#include "kyto_gpu.h"

namespace kg {

// An error inside the library: the status the entry point returns, and its message.
struct Error {
  kg_status status;
  std::string message;
};

[[noreturn]] inline void fail(kg_status status, std::string message) {
  throw Error{status, std::move(message)};
}

[[noreturn]] inline void fail_cuda(cudaError_t e, const char* what, const char* file,
                                   int line) {
  kg_status s = (e == cudaErrorMemoryAllocation) ? KG_ERR_OOM : KG_ERR_DEVICE;
  std::string msg = std::string("CUDA error ") + cudaGetErrorName(e) + " (" +
                    cudaGetErrorString(e) + ") in " + what + " at " + file + ":" +
                    std::to_string(line);
  if (s == KG_ERR_OOM) msg += "; the device ran out of memory: lower memory_limit";
  fail(s, msg);
}

#define KG_CUDA(call)                                                   \
  do {                                                                  \
    cudaError_t kg_e_ = (call);                                         \
    if (kg_e_ != cudaSuccess) ::kg::fail_cuda(kg_e_, #call, __FILE__, __LINE__); \
  } while (0)

#define KG_CUBLAS(call)                                                            \
  do {                                                                             \
    cublasStatus_t kg_s_ = (call);                                                 \
    if (kg_s_ != CUBLAS_STATUS_SUCCESS)                                            \
      ::kg::fail(KG_ERR_DEVICE, std::string("cuBLAS status ") +                    \
                                    std::to_string((int)kg_s_) + " in " #call);    \
  } while (0)

#define KG_CUSOLVER(call)                                                          \
  do {                                                                             \
    cusolverStatus_t kg_s_ = (call);                                               \
    if (kg_s_ != CUSOLVER_STATUS_SUCCESS)                                          \
      ::kg::fail(KG_ERR_DEVICE, std::string("cuSOLVER status ") +                  \
                                    std::to_string((int)kg_s_) + " in " #call);    \
  } while (0)

// Kernels of this library launched so far (kg_diag_kernel_launches); every launch
// site is followed by KG_LAUNCH_CHECK.
extern std::atomic<uint64_t> g_launches;

#define KG_LAUNCH_CHECK()                        \
  do {                                           \
    ::kg::g_launches.fetch_add(1, std::memory_order_relaxed); \
    KG_CUDA(cudaGetLastError());                 \
  } while (0)

// The calling thread's last error message (kg_last_error).
std::string& last_error();

// Whether KYTO_GPU_TRACE is set (read once).
inline bool trace_on() {
  static const bool on = std::getenv("KYTO_GPU_TRACE") != nullptr;
  return on;
}

// Under KYTO_GPU_TRACE, an allocation whose host call took over 2 ms is reported with
// its size and the device pool's reserved and used bytes after it (the pool grows, and
// the call blocks, when no free range of the pool fits the request).
void trace_slow_alloc(size_t bytes, double ms);

// The library's own stream-ordered memory pool on `device` (created at the first use,
// kept until the process ends), with its release threshold at the maximum: memory this
// library frees stays with its pool for the next call instead of going back to the
// driver, and no other allocator's pool (the device's default pool, which a PyTorch or
// CuPy process may use) has its threshold changed.
cudaMemPool_t device_pool(int device);

// Allocation failures injected for tests (kg_diag_fail_allocations): after `n` more
// allocations every allocation fails as out of memory, until the count is reset.
extern std::atomic<uint64_t> g_allocs_left;

// A device allocation, stream-ordered (cudaMallocFromPoolAsync on the library's pool /
// cudaFreeAsync).
template <class T>
struct DeviceBuffer {
  T* ptr = nullptr;
  size_t count = 0;
  cudaStream_t stream = nullptr;

  DeviceBuffer() = default;
  DeviceBuffer(size_t n, cudaStream_t s) { alloc(n, s); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept { swap(o); }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    reset();
    swap(o);
    return *this;
  }
  ~DeviceBuffer() { reset(); }

  void swap(DeviceBuffer& o) noexcept {
    std::swap(ptr, o.ptr);
    std::swap(count, o.count);
    std::swap(stream, o.stream);
  }
  void alloc(size_t n, cudaStream_t s) {
    reset();
    stream = s;
    count = n;
    if (!n) return;
    if (g_allocs_left.load(std::memory_order_relaxed) != UINT64_MAX) {
      uint64_t left = g_allocs_left.load();
      while (left != UINT64_MAX && left > 0 && !g_allocs_left.compare_exchange_weak(left, left - 1)) {
      }
      if (left == 0) {
        count = 0;
        fail_cuda(cudaErrorMemoryAllocation, "an injected allocation failure", __FILE__, __LINE__);
      }
    }
    int device = 0;
    KG_CUDA(cudaGetDevice(&device));
    cudaMemPool_t pool = device_pool(device);
    if (!trace_on()) {
      KG_CUDA(cudaMallocFromPoolAsync((void**)&ptr, n * sizeof(T), pool, s));
      return;
    }
    auto t0 = std::chrono::steady_clock::now();
    KG_CUDA(cudaMallocFromPoolAsync((void**)&ptr, n * sizeof(T), pool, s));
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (ms > 2.0) trace_slow_alloc(n * sizeof(T), ms);
  }
  void reset() noexcept {
    if (ptr) cudaFreeAsync(ptr, stream);
    ptr = nullptr;
    count = 0;
  }
  void zero() {
    if (count) KG_CUDA(cudaMemsetAsync(ptr, 0, count * sizeof(T), stream));
  }
  T* get() const { return ptr; }
  size_t bytes() const { return count * sizeof(T); }
};

// Whether p is memory the device can read directly (device or managed).
inline bool is_device_pointer(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a{};
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Whether p is ordinary (pageable) host memory: neither the device's nor page-locked.
inline bool is_pageable_host(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a{};
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

// Copies `bytes` of pageable host memory to the device through page-locked staging
// buffers of this process (two 16 MB halves, filled by the host while the other half's
// copy runs on `stream`), so that copies from several host threads run side by side at
// the link's rate instead of through the driver's own staging. Returns once every byte
// has been read from `src` and the staging buffers are free again (kg_context.cu).
void staged_copy_to_device(void* dst, const void* src, size_t bytes, cudaStream_t stream);

// Set in the batching form's worker threads: their pageable copies go through the
// staging buffers. A single caller keeps the driver's own pageable copy, which is faster
// than one host thread filling the staging buffers; several workers filling their own
// staging buffers side by side are faster than the driver's copies, which serialize.
extern thread_local bool g_stage_pageable;

// `count` elements at `src` (host or device) as a device pointer: src itself when the
// device can read it, else a copy in `holder` (in a batching worker, pageable sources of
// 4 MB or more through the staging buffers).
template <class T>
const T* device_view(const T* src, size_t count, DeviceBuffer<T>& holder,
                     cudaStream_t stream) {
  if (is_device_pointer(src)) return src;
  holder.alloc(count, stream);
  const size_t bytes = count * sizeof(T);
  if (g_stage_pageable && bytes >= (4u << 20) && is_pageable_host(src))
    staged_copy_to_device(holder.ptr, src, bytes, stream);
  else if (count)
    KG_CUDA(cudaMemcpyAsync(holder.ptr, src, bytes, cudaMemcpyHostToDevice, stream));
  return holder.ptr;
}

}  // namespace kg

// The context behind the C ABI's kg_ctx.
struct kg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cublasHandle_t cublas = nullptr;
  cusolverDnHandle_t cusolver = nullptr;
  std::mutex handles;  // cuBLAS/cuSOLVER handles are bound to one stream at a time
  // Session resources (a stream with its own cuBLAS and cuSOLVER handles) returned by
  // finished PCA sessions, reused by the next: creating and destroying the handles
  // (and their workspaces) costs far more than a session's dense steps.
  struct SessionRes {
    cudaStream_t stream = nullptr;
    cublasHandle_t cublas = nullptr;
    cusolverDnHandle_t cusolver = nullptr;
  };
  std::mutex res_mu;
  std::vector<SessionRes> free_res;
  // The exact kNN's candidate slices (n x 512 keys and rows: 16 GB at 4M rows), kept and
  // grown between calls so a search does not wait on the pool for them; the searches
  // of one context run one at a time on its stream.
  kg::DeviceBuffer<uint8_t> knn_ws;
  const volatile int32_t* cancel = nullptr;
  std::atomic<uint64_t> done{0}, total{0};
  int sm_count = 0;
  // Seconds a bounded wait gives the device before KG_ERR_TIMEOUT.
  double wait_limit_s = 900.0;
};

namespace kg {

// Make ctx's device current for this thread.
inline void use_device(kg_ctx* ctx) { KG_CUDA(cudaSetDevice(ctx->device)); }

inline void check_cancel(const kg_ctx* ctx) {
  if (ctx->cancel && *ctx->cancel) fail(KG_CANCELLED, "the run was cancelled");
}

// Wait for `stream` with a deadline: polls an event instead of blocking forever, so a
// stuck device surfaces as KG_ERR_TIMEOUT, and the cancel flag is honoured meanwhile
// (the work already queued still runs to its end before the call returns).
inline void wait_stream(kg_ctx* ctx, cudaStream_t stream) {
  cudaEvent_t ev;
  KG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  KG_CUDA(cudaEventRecord(ev, stream));
  auto start = std::chrono::steady_clock::now();
  int spins = 0;
  for (;;) {
    cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) {
      cudaEventDestroy(ev);
      fail_cuda(e, "cudaEventQuery (a kernel failed)", __FILE__, __LINE__);
    }
    double waited =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    if (waited > ctx->wait_limit_s) {
      cudaEventDestroy(ev);
      fail(KG_ERR_TIMEOUT, "the device did not finish within the wait limit");
    }
    if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  cudaEventDestroy(ev);
}

// Phase timings of a call, on its stream, printed to stderr when KYTO_GPU_TRACE is set
// (one line per call: phase name, count, device ms between the stream's marks, and the
// host's wall ms between the same marks; a host figure far above the device one means
// the stream sat idle while the host worked or waited). Costs nothing when unset.
struct Trace {
  bool on = false;
  cudaStream_t s = nullptr;
  std::string what;
  struct Mark {
    std::string name;
    cudaEvent_t ev;
    std::chrono::steady_clock::time_point host;
  };
  std::vector<Mark> marks;
  Trace(cudaStream_t st, const char* call) : s(st), what(call) {
    on = trace_on();
    mark("start");
  }
  void mark(const char* name) {
    if (!on) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, s);
    marks.push_back({name, e, std::chrono::steady_clock::now()});
  }
  ~Trace() {
    if (!on || marks.empty()) return;
    cudaEventSynchronize(marks.back().ev);
    struct Acc {
      std::string name;
      int n;
      double dev, host;
    };
    std::vector<Acc> acc;
    for (size_t i = 1; i < marks.size(); ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, marks[i - 1].ev, marks[i].ev);
      double host =
          std::chrono::duration<double, std::milli>(marks[i].host - marks[i - 1].host).count();
      bool found = false;
      for (auto& a : acc)
        if (a.name == marks[i].name) {
          a.n += 1;
          a.dev += ms;
          a.host += host;
          found = true;
        }
      if (!found) acc.push_back({marks[i].name, 1, ms, host});
    }
    std::string line = "[kyto_gpu trace] " + what + ":";
    for (auto& a : acc) {
      char buf[160];
      std::snprintf(buf, sizeof buf, " %s x%d %.3f ms (host %.3f);", a.name.c_str(), a.n, a.dev,
                    a.host);
      line += buf;
    }
    std::fprintf(stderr, "%s\n", line.c_str());
    for (auto& m : marks) cudaEventDestroy(m.ev);
  }
};

template <class F>
kg_status guarded(F&& body) {
  try {
    body();
    return KG_OK;
  } catch (const Error& e) {
    last_error() = e.message;
    return e.status;
  } catch (const std::bad_alloc&) {
    last_error() = "host memory exhausted";
    return KG_ERR_OOM;
  } catch (const std::exception& e) {
    last_error() = e.what();
    return KG_ERR_DEVICE;
  } catch (...) {
    last_error() = "unknown error";
    return KG_ERR_DEVICE;
  }
}

inline unsigned blocks_for(uint64_t n, unsigned per_block) {
  uint64_t b = (n + per_block - 1) / per_block;
  return (unsigned)(b ? b : 1);
}

}  // namespace kg
