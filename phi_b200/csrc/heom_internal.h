// heom_internal.h -- host-side internals shared by the library's translation
// units (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "heom_device.cuh"

namespace phi {

// Device / pinned host allocations reused across contexts of the process
// (device_cache.cpp).
cudaError_t cached_device_alloc(void **out, size_t bytes);
void cached_device_free(void *p, size_t bytes);
cudaError_t cached_host_alloc(void **out, size_t bytes);
void cached_host_free(void *p, size_t bytes);

// Owning device allocation (through the process-level cache).
struct DeviceBuffer {
  void *ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&o) noexcept : ptr(o.ptr), bytes(o.bytes) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
    if (this != &o) {
      reset();
      ptr = o.ptr;
      bytes = o.bytes;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DeviceBuffer() { reset(); }
  cudaError_t alloc(size_t n) {
    reset();
    if (n == 0) n = 16;
    cudaError_t e = cached_device_alloc(&ptr, n);
    if (e != cudaSuccess) {
      ptr = nullptr;
      return e;
    }
    bytes = n;
    return cudaSuccess;
  }
  void reset() {
    if (ptr) cached_device_free(ptr, bytes);
    ptr = nullptr;
    bytes = 0;
  }
  template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Result of the device hierarchy construction.
struct DeviceHierarchy {
  int64_t M = 0;
  int T = 0;
  int L = 0;
  int64_t budget = 0;  // node budget; 0 = none
  std::vector<long long> tier_count;
  std::vector<long long> tier_first;
  DeviceBuffer mi;          // M*T uint8
  DeviceBuffer next;        // M*T int32
  DeviceBuffer prev;        // M*T int32
  DeviceBuffer rank_to_id;  // M int32, per tier by colex rank
};

// Builds PHI's node order and neighbour tables on the device.  Returns 0 or a
// PHI_E_* style code (2 = OOM, 3 = budget, 7 = CUDA, 1 = invalid).
int build_hierarchy_device(int T, int L, DeviceHierarchy *out, std::string *err,
                           cudaStream_t stream);

}  // namespace phi
