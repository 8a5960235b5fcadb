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

struct DevArena {
  std::vector<void *> ptrs;
  long long bytes = 0;
  cudaError_t err = cudaSuccess;
  // zero-filled unless the caller overwrites it at once (upload)
  template <typename T>
  T *alloc(size_t count, bool zero = true) {
    if (count == 0) count = 1;
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      err = e;
      return nullptr;
    }
    if (zero) cudaMemset(p, 0, count * sizeof(T));
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
    for (void *p : ptrs) cudaFree(p);
    ptrs.clear();
    bytes = 0;
  }
  ~DevArena() { release(); }
};

}  // namespace clgpu
