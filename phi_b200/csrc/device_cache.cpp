// device_cache.cpp -- reuse of device (and small pinned host) allocations
// across contexts in one process.
//
// A user job that builds a context, propagates and destroys it pays a dozen
// or more cudaMalloc / cudaFree pairs; on a shared machine each of those can
// take milliseconds.  Freed blocks are kept per (device, size) and handed to
// the next allocation of exactly that size, as a caching allocator does.  A
// free still synchronises the device first (the guarantee cudaFree gives),
// so no block is reused while a kernel of its previous owner runs; blocks
// are filed under the device they live on.  At most
// kMaxCachedBytes stay cached; an allocation that fails with out-of-memory
// releases the cache and retries; phi_gpu_release_cached_memory releases it
// on request.  Nothing is released at process exit (the driver reclaims it).
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/phi_b200.h"
#include "heom_internal.h"

namespace phi {
namespace {

constexpr size_t kMaxCachedBytes = size_t(8) << 30;

struct Cache {
  std::mutex mu;
  std::map<std::pair<int, size_t>, std::vector<void *>> dev;  // (device, bytes) -> blocks
  std::map<size_t, std::vector<void *>> host;                  // pinned host blocks by size
  size_t dev_bytes = 0;
};

Cache &cache() {
  static Cache *c = new Cache();  // never destroyed: frees at exit would race the runtime
  return *c;
}

size_t release_device_locked(Cache &c, int device) {
  size_t freed = 0;
  for (auto it = c.dev.begin(); it != c.dev.end();) {
    if (device >= 0 && it->first.first != device) {
      ++it;
      continue;
    }
    for (void *p : it->second) {
      cudaFree(p);
      freed += it->first.second;
    }
    c.dev_bytes -= it->first.second * it->second.size();
    it = c.dev.erase(it);
  }
  return freed;
}

}  // namespace

cudaError_t cached_device_alloc(void **out, size_t bytes) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  Cache &c = cache();
  {
    std::lock_guard<std::mutex> lock(c.mu);
    auto it = c.dev.find({device, bytes});
    if (it != c.dev.end() && !it->second.empty()) {
      *out = it->second.back();
      it->second.pop_back();
      c.dev_bytes -= bytes;
      return cudaSuccess;
    }
  }
  e = cudaMalloc(out, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // clear the recorded error before the retry
    {
      std::lock_guard<std::mutex> lock(c.mu);
      release_device_locked(c, device);
    }
    e = cudaMalloc(out, bytes);
  }
  return e;
}

void cached_device_free(void *p, size_t bytes) {
  if (!p) return;
  // The block is filed under the device it lives on (the current device may
  // have changed since it was allocated), after that device has finished
  // its work.
  cudaPointerAttributes attr{};
  int current = 0;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess || attr.type != cudaMemoryTypeDevice ||
      cudaGetDevice(&current) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(p);
    return;
  }
  const int device = attr.device;
  bool synced = true;
  if (device != current) synced = cudaSetDevice(device) == cudaSuccess;
  synced = synced && cudaDeviceSynchronize() == cudaSuccess;
  if (device != current) cudaSetDevice(current);
  if (!synced) {
    cudaFree(p);
    return;
  }
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  if (c.dev_bytes + bytes > kMaxCachedBytes) {
    cudaFree(p);
    return;
  }
  c.dev[{device, bytes}].push_back(p);
  c.dev_bytes += bytes;
}

cudaError_t cached_host_alloc(void **out, size_t bytes) {
  Cache &c = cache();
  {
    std::lock_guard<std::mutex> lock(c.mu);
    auto it = c.host.find(bytes);
    if (it != c.host.end() && !it->second.empty()) {
      *out = it->second.back();
      it->second.pop_back();
      return cudaSuccess;
    }
  }
  return cudaMallocHost(out, bytes);
}

void cached_host_free(void *p, size_t bytes) {
  if (!p) return;
  Cache &c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  auto &v = c.host[bytes];
  if (v.size() >= 64) {
    cudaFreeHost(p);
    return;
  }
  v.push_back(p);
}

}  // namespace phi

extern "C" int64_t phi_gpu_release_cached_memory(void) {
  phi::Cache &c = phi::cache();
  std::lock_guard<std::mutex> lock(c.mu);
  const size_t freed = phi::release_device_locked(c, -1);
  for (auto &kv : c.host)
    for (void *p : kv.second) cudaFreeHost(p);
  c.host.clear();
  return (int64_t)freed;
}
