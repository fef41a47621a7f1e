// Caching allocator for handle arenas, batch tables and pinned control blocks.
#include "alloc.h"

#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/fluid_pp.h"

namespace fpp {
void set_global_error(const std::string& message);
}

namespace {

constexpr int kHostKey = -1;   // cache key of pinned host memory

struct Cache {
  size_t limit = 0;     // bytes the free list may hold (0: caching off)
  size_t cached = 0;    // bytes on the free list
  std::multimap<size_t, void*> blocks;   // free blocks by size
};

struct Live {
  int key;
  size_t bytes;
};

std::mutex g_mu;
std::map<int, Cache> g_cache;
std::unordered_map<void*, Live> g_live;

// Block sizes: powers of two up to 1 MiB, then multiples of 2 MiB, so that
// handles of nearby sizes share blocks.
size_t block_size(size_t bytes) {
  constexpr size_t kSmall = size_t(1) << 20, kGrain = size_t(2) << 20;
  if (bytes <= kSmall) {
    size_t s = 256;
    while (s < bytes) s <<= 1;
    return s;
  }
  return (bytes + kGrain - 1) / kGrain * kGrain;
}

void raw_free(int key, void* p) {
  if (key == kHostKey) cudaFreeHost(p);
  else cudaFree(p);
}

cudaError_t raw_alloc(int key, void** p, size_t bytes) {
  return key == kHostKey ? cudaMallocHost(p, bytes) : cudaMalloc(p, bytes);
}

// Frees the free list of `key` down to `keep` bytes (caller holds no lock).
void trim(int key, size_t keep) {
  std::vector<void*> out;
  {
    std::lock_guard<std::mutex> g(g_mu);
    Cache& c = g_cache[key];
    while (c.cached > keep && !c.blocks.empty()) {
      auto it = std::prev(c.blocks.end());   // largest first
      c.cached -= it->first;
      out.push_back(it->second);
      c.blocks.erase(it);
    }
  }
  for (void* p : out) raw_free(key, p);
}

cudaError_t alloc_key(int key, void** p, size_t bytes) {
  const size_t bs = block_size(bytes ? bytes : 1);
  {
    std::lock_guard<std::mutex> g(g_mu);
    Cache& c = g_cache[key];
    auto it = c.blocks.lower_bound(bs);
    if (it != c.blocks.end() && it->first <= bs + bs / 4) {
      *p = it->second;
      g_live[*p] = Live{key, it->first};
      c.cached -= it->first;
      c.blocks.erase(it);
      return cudaSuccess;
    }
  }
  cudaError_t e = raw_alloc(key, p, bs);
  if (e == cudaErrorMemoryAllocation) {   // cached blocks of other sizes may be what is missing
    cudaGetLastError();
    trim(key, 0);
    e = raw_alloc(key, p, bs);
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  std::lock_guard<std::mutex> g(g_mu);
  g_live[*p] = Live{key, bs};
  return cudaSuccess;
}

void release_key(void* p, cudaStream_t last_use) {
  if (!p) return;
  Live info{};
  bool keep = false;
  {
    std::lock_guard<std::mutex> g(g_mu);
    auto it = g_live.find(p);
    if (it == g_live.end()) return;   // not ours
    info = it->second;
    g_live.erase(it);
    const Cache& c = g_cache[info.key];
    keep = c.cached + info.bytes <= c.limit;
  }
  if (!keep) {
    raw_free(info.key, p);
    return;
  }
  cudaStreamSynchronize(last_use);   // the block's last work has finished before anyone reuses it
  std::lock_guard<std::mutex> g(g_mu);
  Cache& c = g_cache[info.key];
  c.blocks.emplace(info.bytes, p);
  c.cached += info.bytes;
}

int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

}  // namespace

namespace fpp {

cudaError_t dev_alloc(void** p, size_t bytes) { return alloc_key(current_device(), p, bytes); }
void dev_release(void* p, cudaStream_t last_use) { release_key(p, last_use); }
cudaError_t host_alloc(void** p, size_t bytes) { return alloc_key(kHostKey, p, bytes); }
void host_release(void* p, cudaStream_t last_use) { release_key(p, last_use); }

}  // namespace fpp

// ------------------------------------------------------------------ C ABI
extern "C" {

int fluid_pp_set_allocation_cache(int device, unsigned long long max_cached_bytes) {
  if (device < kHostKey) return FLUID_PP_INVALID_ARG;
  int prev = 0;
  if (device >= 0) {
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) {
      cudaGetLastError();
      fpp::set_global_error("allocation cache: no such device");
      return FLUID_PP_INVALID_ARG;
    }
  }
  {
    std::lock_guard<std::mutex> g(g_mu);
    g_cache[device].limit = size_t(max_cached_bytes);
  }
  trim(device, size_t(max_cached_bytes));
  if (device >= 0) cudaSetDevice(prev);
  return FLUID_PP_OK;
}

int fluid_pp_allocation_cache_bytes(int device, unsigned long long* cached_bytes) {
  if (device < kHostKey || !cached_bytes) return FLUID_PP_INVALID_ARG;
  std::lock_guard<std::mutex> g(g_mu);
  auto it = g_cache.find(device);
  *cached_bytes = it == g_cache.end() ? 0ull : (unsigned long long)it->second.cached;
  return FLUID_PP_OK;
}

}  // extern "C"
