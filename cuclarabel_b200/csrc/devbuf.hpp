// devbuf.hpp -- owning list of device allocations made at setup time.
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <utility>
#include <vector>

#include "pinned.hpp"

namespace clgpu {

// Host vector of a large setup array: page-locked pool memory, elements
// default-initialised (PinnedInitAlloc).
template <class T>
using hvec = std::vector<T, PinnedInitAlloc<T>>;

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
  bool pending = false;  // uploads not yet settled
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
  // Uploads are asynchronous on the legacy stream, so they overlap the
  // host work that follows.  A page-locked source (an hvec) is copied from
  // in place and kept out of the pool until settle(); a small pageable
  // source is first copied into a page-locked pool buffer (a pageable copy
  // would wait for every copy before it); a large one is copied directly
  // (the call returns once the driver has staged it).  The caller must not
  // change an hvec after uploading it, and must call settle() once it has
  // synchronised the legacy stream.
  template <typename T, typename Al>
  T *upload(const std::vector<T, Al> &v) {
    T *p = alloc<T>(v.size(), v.empty());
    if (p && !v.empty()) copy_in(p, v.data(), v.size() * sizeof(T));
    return p;
  }
  void copy_in(void *dst, const void *src, size_t bytes) {
    constexpr size_t kStageMax = 8u << 20;
    PinnedPool &pool = PinnedPool::get();
    const void *from = src;
    if (pool.owns(src)) {
      pool.hold_for(const_cast<void *>(src), this);
    } else if (bytes <= kStageMax) {
      void *stage = pool.take(bytes);
      if (stage) {
        std::memcpy(stage, src, bytes);
        pool.hold_for(stage, this);
        pool.give(stage);  // returns to the pool at settle()
        from = stage;
      }
    }
    cudaError_t e = cudaMemcpyAsync(dst, from, bytes, cudaMemcpyHostToDevice, 0);
    if (e != cudaSuccess) err = e;
    pending = true;
  }
  // the legacy stream has been synchronised: the upload sources go back
  void settle() {
    PinnedPool::get().settle(this);
    pending = false;
  }
  void release() {
    if (pending) {
      cudaStreamSynchronize(0);
      settle();
    }
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
