// devbuf.hpp -- owning list of device allocations made at setup time.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace clgpu {

struct DevArena {
  std::vector<void *> ptrs;
  long long bytes = 0;
  cudaError_t err = cudaSuccess;
  template <typename T>
  T *alloc(size_t count) {
    if (count == 0) count = 1;
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      err = e;
      return nullptr;
    }
    cudaMemset(p, 0, count * sizeof(T));
    ptrs.push_back(p);
    bytes += (long long)(count * sizeof(T));
    return static_cast<T *>(p);
  }
  template <typename T>
  T *upload(const std::vector<T> &v) {
    T *p = alloc<T>(v.size());
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
