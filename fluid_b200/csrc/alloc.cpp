// Caching allocator for handle arenas, batch tables and pinned control blocks.
//
// Two tiers per device, both used only while caching is on for the device:
//  * slabs reserved up front (fluid_pp_reserve_allocation): device memory
//    handed out by best fit over free address ranges that coalesce on release,
//    so an admission never maps new memory;
//  * a free list of whole blocks from earlier cudaMalloc calls, reused for
//    requests of a similar size (at most a quarter larger).
// Anything else is a plain cudaMalloc / cudaFree.
#include "alloc.h"

#include <iterator>
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

constexpr int kHostKey = -1;     // cache key of pinned host memory
constexpr size_t kAlign = 256;   // slab ranges keep cudaMalloc's alignment

struct Cache {
  size_t limit = 0;     // bytes the block free list may hold (0: caching off)
  size_t cached = 0;    // bytes on the block free list
  std::multimap<size_t, void*> blocks;   // free whole blocks by size
  // slab tier
  std::vector<std::pair<char*, size_t>> slabs;
  std::map<char*, size_t> free_by_addr;        // free ranges by start
  std::multimap<size_t, char*> free_by_size;   // the same ranges by size
};

struct Live {
  int key;
  size_t bytes;
  bool slab;
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

// Slab ranges (caller holds g_mu).
void slab_insert(Cache& c, char* p, size_t n) {
  c.free_by_addr[p] = n;
  c.free_by_size.emplace(n, p);
}
void slab_erase(Cache& c, std::map<char*, size_t>::iterator it) {
  auto range = c.free_by_size.equal_range(it->second);
  for (auto s = range.first; s != range.second; ++s)
    if (s->second == it->first) {
      c.free_by_size.erase(s);
      break;
    }
  c.free_by_addr.erase(it);
}
char* slab_take(Cache& c, size_t n) {
  auto it = c.free_by_size.lower_bound(n);
  if (it == c.free_by_size.end()) return nullptr;
  char* p = it->second;
  const size_t have = it->first;
  slab_erase(c, c.free_by_addr.find(p));
  if (have > n) slab_insert(c, p + n, have - n);
  return p;
}
void slab_give(Cache& c, char* p, size_t n) {
  auto next = c.free_by_addr.lower_bound(p);
  if (next != c.free_by_addr.end() && p + n == next->first) {   // merge with the range after
    n += next->second;
    slab_erase(c, next);
  }
  auto prev = c.free_by_addr.lower_bound(p);
  if (prev != c.free_by_addr.begin()) {
    --prev;
    if (prev->first + prev->second == p) {   // merge with the range before
      p = prev->first;
      n += prev->second;
      slab_erase(c, prev);
    }
  }
  slab_insert(c, p, n);
}

// Frees the block free list of `key` down to `keep` bytes (caller holds no lock).
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
    if (c.limit > 0 && !c.free_by_size.empty()) {
      const size_t n = bytes ? (bytes + kAlign - 1) / kAlign * kAlign : kAlign;
      if (char* s = slab_take(c, n)) {
        *p = s;
        g_live[*p] = Live{key, n, true};
        return cudaSuccess;
      }
    }
    auto it = c.blocks.lower_bound(bs);
    if (it != c.blocks.end() && it->first <= bs + bs / 4) {
      *p = it->second;
      g_live[*p] = Live{key, it->first, false};
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
  g_live[*p] = Live{key, bs, false};
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
    keep = info.slab || c.cached + info.bytes <= c.limit;
  }
  if (!keep) {
    raw_free(info.key, p);
    return;
  }
  cudaStreamSynchronize(last_use);   // the block's last work has finished before anyone reuses it
  std::lock_guard<std::mutex> g(g_mu);
  Cache& c = g_cache[info.key];
  if (info.slab) {
    slab_give(c, static_cast<char*>(p), info.bytes);
  } else {
    c.blocks.emplace(info.bytes, p);
    c.cached += info.bytes;
  }
}

int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

}  // namespace

namespace fpp {

cudaError_t order_streams(cudaStream_t prev, cudaStream_t next) {
  if (prev == next) return cudaSuccess;
  cudaEvent_t ev;
  cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (e != cudaSuccess) return e;
  e = cudaEventRecord(ev, prev);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(next, ev, 0);
  cudaEventDestroy(ev);   // released once the wait has been satisfied
  return e;
}

}  // namespace fpp

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
  std::vector<char*> slabs;
  {
    std::lock_guard<std::mutex> g(g_mu);
    Cache& c = g_cache[device];
    c.limit = size_t(max_cached_bytes);
    // with caching off, the slabs go once none of their ranges is in use
    if (max_cached_bytes == 0) {
      size_t free_bytes = 0, slab_bytes = 0;
      for (const auto& r : c.free_by_addr) free_bytes += r.second;
      for (const auto& s : c.slabs) slab_bytes += s.second;
      if (free_bytes == slab_bytes) {
        for (const auto& s : c.slabs) slabs.push_back(s.first);
        c.slabs.clear();
        c.free_by_addr.clear();
        c.free_by_size.clear();
      }
    }
  }
  trim(device, size_t(max_cached_bytes));
  for (char* s : slabs) raw_free(device, s);
  if (device >= 0) cudaSetDevice(prev);
  return FLUID_PP_OK;
}

int fluid_pp_reserve_allocation(int device, unsigned long long bytes) {
  if (device < 0 || bytes == 0) return FLUID_PP_INVALID_ARG;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    fpp::set_global_error("reserve allocation: no such device");
    return FLUID_PP_INVALID_ARG;
  }
  void* p = nullptr;
  const size_t n = (size_t(bytes) + kAlign - 1) / kAlign * kAlign;
  const cudaError_t e = cudaMalloc(&p, n);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    fpp::set_global_error(std::string("reserve allocation: ") + cudaGetErrorString(e));
    return FLUID_PP_OOM;
  }
  std::lock_guard<std::mutex> g(g_mu);
  Cache& c = g_cache[device];
  c.slabs.emplace_back(static_cast<char*>(p), n);
  slab_give(c, static_cast<char*>(p), n);
  return FLUID_PP_OK;
}

int fluid_pp_allocation_cache_bytes(int device, unsigned long long* cached_bytes) {
  if (device < kHostKey || !cached_bytes) return FLUID_PP_INVALID_ARG;
  std::lock_guard<std::mutex> g(g_mu);
  auto it = g_cache.find(device);
  size_t n = 0;
  if (it != g_cache.end()) {
    n = it->second.cached;
    for (const auto& r : it->second.free_by_addr) n += r.second;
  }
  *cached_bytes = (unsigned long long)n;
  return FLUID_PP_OK;
}

}  // extern "C"
