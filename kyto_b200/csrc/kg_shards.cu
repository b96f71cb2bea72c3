// The shards of kyto's tiled layers decoded on the host, straight into the buffers the
// tile join reads (page-locked ones for the device copies that follow): the read side
// of the Zarr v3 `sharding_indexed` codec with zstd inner chunks that kyto's store uses
// for a layer's indptr, indices and data (docs/format.md 4.4), and the plain
// [bytes, zstd] chunks of tile_offsets. kyto reads them through a third-party Zarr crate;
// this file restates the published layout. Host code only: no kernel.
//
// A shard: its inner chunks' zstd frames back to back, then the index: one
// (offset, nbytes) pair of little-endian u64 per inner chunk in chunk order (both
// 2^64 - 1 for a chunk that is not stored: it reads as the fill value 0), then the
// CRC-32C of the index bytes (little-endian u32). Every inner chunk decodes to the full
// chunk shape (Zarr's regular grid pads the edges with the fill value).
//
// The chunks of one read decode on several host threads (one chunk at a time each,
// handed out in chunk order): KYTO_GPU_DECODE_THREADS, else every hardware thread, for
// reads of 4 MB or more. A failing chunk stops the hand-out; the chunks already handed
// out finish, so the lowest failing chunk is always found and reported, the same on
// every run.
//
// zstd comes from the system's libzstd.so.1, loaded at the first decode (dlopen), so the
// library itself links no compression code and loads where libzstd is absent; a decode
// then fails with KG_ERR_STORE naming the missing library.

#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "kg_internal.cuh"

namespace kg {
namespace {

constexpr uint64_t kMissing = ~0ull;

// CRC-32C (Castagnoli): reflected polynomial 0x82F63B78, initial and final XOR all ones.
struct Crc32cTable {
  uint32_t t[256];
  constexpr Crc32cTable() : t{} {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1u) ? (c >> 1) ^ 0x82F63B78u : c >> 1;
      t[i] = c;
    }
  }
};
constexpr Crc32cTable kCrc32c{};

uint32_t crc32c(const uint8_t* p, size_t n) {
  uint32_t c = 0xFFFFFFFFu;
  for (size_t i = 0; i < n; ++i) c = kCrc32c.t[(c ^ p[i]) & 0xFFu] ^ (c >> 8);
  return c ^ 0xFFFFFFFFu;
}

uint64_t le64(const uint8_t* p) {
  uint64_t v = 0;
  for (int i = 7; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}

uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// libzstd's one-shot decoder, looked up once.
struct Zstd {
  size_t (*decompress)(void*, size_t, const void*, size_t) = nullptr;
  unsigned (*is_error)(size_t) = nullptr;
  const char* (*error_name)(size_t) = nullptr;
  std::string why;
};

const Zstd& zstd() {
  static const Zstd z = [] {
    Zstd z;
    void* h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
      const char* e = dlerror();
      z.why = std::string("libzstd.so.1 could not be loaded (") + (e ? e : "?") + ")";
      return z;
    }
    z.decompress = reinterpret_cast<size_t (*)(void*, size_t, const void*, size_t)>(
        dlsym(h, "ZSTD_decompress"));
    z.is_error = reinterpret_cast<unsigned (*)(size_t)>(dlsym(h, "ZSTD_isError"));
    z.error_name = reinterpret_cast<const char* (*)(size_t)>(dlsym(h, "ZSTD_getErrorName"));
    if (!z.decompress || !z.is_error || !z.error_name) {
      z.decompress = nullptr;
      z.why = "libzstd.so.1 lacks ZSTD_decompress";
    }
    return z;
  }();
  return z;
}

[[noreturn]] void store_fail(const std::string& detail) {
  fail(KG_ERR_STORE, "could not read the shard: " + detail);
}

// One zstd frame that must decode to exactly `bytes` bytes.
void decode_frame(const uint8_t* src, size_t n, void* dst, size_t bytes, uint64_t chunk) {
  const Zstd& z = zstd();
  if (!z.decompress) store_fail(z.why);
  const size_t got = z.decompress(dst, bytes, src, n);
  if (z.is_error(got))
    store_fail("inner chunk " + std::to_string(chunk) + ": zstd: " + z.error_name(got));
  if (got != bytes)
    store_fail("inner chunk " + std::to_string(chunk) + " decodes to " + std::to_string(got) +
               " bytes, not the chunk's " + std::to_string(bytes));
}

}  // namespace
}  // namespace kg

using namespace kg;

extern "C" {

kg_status kg_shard_read(const uint8_t* shard, uint64_t shard_bytes, uint64_t chunks_per_shard,
                        uint64_t chunk_elems, uint32_t elem_bytes, uint64_t first,
                        uint64_t count, void* out) {
  return guarded([&] {
    if ((!shard && shard_bytes) || (!out && count))
      fail(KG_ERR_INVALID, "kg_shard_read: NULL argument");
    if (elem_bytes != 4 && elem_bytes != 8)
      fail(KG_ERR_INVALID, "kg_shard_read: elements of 4 or 8 bytes");
    if (chunk_elems == 0 || chunks_per_shard == 0 || chunks_per_shard > (1ull << 40))
      fail(KG_ERR_INVALID, "kg_shard_read: a shard of at least one chunk of one element");
    const unsigned __int128 span = (unsigned __int128)chunks_per_shard * chunk_elems;
    if ((unsigned __int128)first + count > span)
      fail(KG_ERR_INVALID, "kg_shard_read: elements past the shard's " +
                               std::to_string((uint64_t)span));
    if ((unsigned __int128)chunk_elems * elem_bytes > (1ull << 40))
      fail(KG_ERR_INVALID, "kg_shard_read: an inner chunk above 2^40 bytes");
    const uint64_t index_bytes = 16 * chunks_per_shard + 4;
    if (shard_bytes < index_bytes)
      store_fail("it holds " + std::to_string(shard_bytes) + " bytes, fewer than its index's " +
                 std::to_string(index_bytes));
    const uint64_t body = shard_bytes - index_bytes;
    const uint8_t* index = shard + body;
    if (crc32c(index, 16 * chunks_per_shard) != le32(index + 16 * chunks_per_shard))
      store_fail("the index's CRC-32C does not match");
    if (!count) return;
    const uint64_t chunk_bytes = chunk_elems * elem_bytes;
    uint8_t* dst = static_cast<uint8_t*>(out);
    const uint64_t last = first + count - 1;
    const uint64_t c_first = first / chunk_elems, c_last = last / chunk_elems;
    // One chunk: its elements that the range holds, decoded into their place in `out`.
    auto one = [&](uint64_t c, std::vector<uint8_t>& scratch) {
      const uint64_t off = le64(index + 16 * c), nb = le64(index + 16 * c + 8);
      const uint64_t lo = std::max(first, c * chunk_elems);
      const uint64_t hi = std::min(last + 1, (c + 1) * chunk_elems);
      uint8_t* to = dst + (lo - first) * elem_bytes;
      if (off == kMissing && nb == kMissing) {
        std::memset(to, 0, (hi - lo) * elem_bytes);
        return;
      }
      if (off == kMissing || nb == kMissing || off > body || nb > body - off)
        store_fail("inner chunk " + std::to_string(c) + " lies outside the shard's " +
                   std::to_string(body) + " bytes of chunks");
      if (lo == c * chunk_elems && hi == (c + 1) * chunk_elems) {
        decode_frame(shard + off, nb, to, chunk_bytes, c);  // the whole chunk, in place
      } else {
        scratch.resize(chunk_bytes);
        decode_frame(shard + off, nb, scratch.data(), chunk_bytes, c);
        std::memcpy(to, scratch.data() + (lo - c * chunk_elems) * elem_bytes,
                    (hi - lo) * elem_bytes);
      }
    };
    const uint64_t n_chunks = c_last - c_first + 1;
    unsigned threads = std::max(1u, std::thread::hardware_concurrency());
    if (const char* t = std::getenv("KYTO_GPU_DECODE_THREADS")) threads = std::max(1, std::atoi(t));
    if (count * elem_bytes < (4u << 20)) threads = 1;
    threads = (unsigned)std::min<uint64_t>(threads, n_chunks);
    std::atomic<uint64_t> next{c_first};
    std::atomic<bool> stop{false};
    // Per thread: the lowest chunk that failed on it and the error.
    std::vector<uint64_t> bad(threads, kMissing);
    std::vector<Error> errors(threads);
    auto work = [&](unsigned t) {
      std::vector<uint8_t> scratch;
      while (!stop.load(std::memory_order_relaxed)) {
        const uint64_t c = next.fetch_add(1);
        if (c > c_last) break;
        // Nothing may leave a worker: an exception escaping a thread ends the process.
        Error err;
        bool failed = true;
        try {
          one(c, scratch);
          failed = false;
        } catch (const Error& e) {
          err = e;
        } catch (const std::bad_alloc&) {
          err = Error{KG_ERR_OOM, "host memory exhausted while decoding inner chunk " +
                                      std::to_string(c)};
        } catch (...) {
          err = Error{KG_ERR_STORE, "could not read the shard: inner chunk " +
                                        std::to_string(c) + ": an unknown error"};
        }
        if (failed) {
          if (c < bad[t]) {
            bad[t] = c;
            errors[t] = err;
          }
          stop.store(true);
        }
      }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < threads; ++t) {
      // A thread that cannot be started leaves its chunks to the others (the calling
      // thread takes part in the hand-out too), never a joinable thread behind a throw.
      try {
        pool.emplace_back(work, t);
      } catch (...) {
        break;
      }
    }
    work(0);
    for (auto& th : pool) th.join();
    unsigned worst = 0;
    for (unsigned t = 1; t < threads; ++t)
      if (bad[t] < bad[worst]) worst = t;
    if (bad[worst] != kMissing) throw errors[worst];
  });
}

kg_status kg_chunk_read(const uint8_t* chunk, uint64_t chunk_bytes, uint64_t elems,
                        uint32_t elem_bytes, void* out) {
  return guarded([&] {
    if (!chunk || !out) fail(KG_ERR_INVALID, "kg_chunk_read: NULL argument");
    if (elem_bytes != 4 && elem_bytes != 8)
      fail(KG_ERR_INVALID, "kg_chunk_read: elements of 4 or 8 bytes");
    if (elems == 0 || (unsigned __int128)elems * elem_bytes > (1ull << 40))
      fail(KG_ERR_INVALID, "kg_chunk_read: a chunk of 1 element to 2^40 bytes");
    decode_frame(chunk, chunk_bytes, out, elems * elem_bytes, 0);
  });
}

}  // extern "C"
