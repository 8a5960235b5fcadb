// devbuf.hpp -- owning list of device allocations made at setup time.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <utility>
#include <vector>

namespace clgpu {

// Host vector whose elements are default-initialised (no zero fill): large
// setup arrays are written in full by parallel threads, so the zeroing pass
// (serial, and the first touch of every page) is skipped.
template <class T>
struct DefaultInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = DefaultInitAlloc<U>;
  };
  DefaultInitAlloc() = default;
  template <class U>
  DefaultInitAlloc(const DefaultInitAlloc<U> &) {}
  template <class U>
  void construct(U *p) noexcept {
    ::new (static_cast<void *>(p)) U;
  }
  template <class U, class... Args>
  void construct(U *p, Args &&...args) {
    ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
  }
};
template <class T>
using hvec = std::vector<T, DefaultInitAlloc<T>>;

// Where the device has memory pools, allocations come from the
// stream-ordered pool on the legacy stream (cudaMallocAsync) and go back
// with cudaFreeAsync, which does not synchronise the device: a solver can
// be set up and destroyed while other solvers run on their own streams
// (serving).  The owner must have no work of its own pending on another
// stream when it releases (every solver entry point that launches work
// finishes it or leaves it to a stream the caller synchronises before
// destroying).  Plain cudaMalloc / cudaFree otherwise.
inline bool arena_pool_alloc() {
  static const bool on = [] {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMemoryPoolsSupported, dev) != cudaSuccess)
      return false;
    if (v == 0) return false;
    // keep freed memory in the pool (no unmapping at each synchronisation;
    // solvers set up and destroyed while others run reuse it)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      unsigned long long keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    return true;
  }();
  return on;
}

struct DevArena {
  std::vector<void *> ptrs;
  long long bytes = 0;
  cudaError_t err = cudaSuccess;
  bool pooled = arena_pool_alloc();
  // zero-filled unless the caller overwrites it at once (upload); ordered
  // on the legacy stream, which the setup synchronises before returning
  template <typename T>
  T *alloc(size_t count, bool zero = true) {
    if (count == 0) count = 1;
    void *p = nullptr;
    cudaError_t e = pooled ? cudaMallocAsync(&p, count * sizeof(T), 0)
                           : cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      err = e;
      return nullptr;
    }
    if (zero) cudaMemsetAsync(p, 0, count * sizeof(T), 0);
    ptrs.push_back(p);
    bytes += (long long)(count * sizeof(T));
    return static_cast<T *>(p);
  }
  template <typename T, typename Al>
  T *upload(const std::vector<T, Al> &v) {
    T *p = alloc<T>(v.size(), v.empty());
    if (p && !v.empty()) {
      cudaError_t e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) err = e;
    }
    return p;
  }
  void release() {
    for (void *p : ptrs) {
      if (pooled)
        cudaFreeAsync(p, 0);
      else
        cudaFree(p);
    }
    ptrs.clear();
    bytes = 0;
  }
  ~DevArena() { release(); }
};

}  // namespace clgpu
