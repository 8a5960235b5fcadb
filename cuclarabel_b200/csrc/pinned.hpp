// pinned.hpp -- page-locked host buffers from a process-wide pool.
//
// cudaFreeHost synchronises the whole device, so a solver destroyed while
// others run on their own streams (serving: a cohort freed while the
// resident lanes step) would stall every stream until the device is idle.
// Buffers released here go back to a pool keyed by their size class (powers
// of two from 256 bytes) and are reused by later solvers; the pool keeps
// its memory for the life of the process.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <map>
#include <mutex>
#include <vector>

namespace clgpu {

class PinnedPool {
 public:
  static PinnedPool &get() {
    static PinnedPool *p = new PinnedPool();  // never destroyed: no cudaFreeHost at exit
    return *p;
  }
  // a buffer of at least `bytes` bytes, or nullptr when the allocation fails
  void *take(size_t bytes) {
    const size_t cls = size_class(bytes);
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto &fl = free_[cls];
      if (!fl.empty()) {
        void *p = fl.back();
        fl.pop_back();
        cls_of_[p] = cls;
        return p;
      }
    }
    void *p = nullptr;
    if (cudaMallocHost(&p, cls) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu_);
    cls_of_[p] = cls;
    return p;
  }
  void give(void *p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu_);
    auto it = cls_of_.find(p);
    if (it == cls_of_.end()) return;
    free_[it->second].push_back(p);
    cls_of_.erase(it);
  }

 private:
  static size_t size_class(size_t bytes) {
    size_t c = 256;
    while (c < bytes) c <<= 1;
    return c;
  }
  std::mutex mu_;
  std::map<size_t, std::vector<void *>> free_;
  std::map<void *, size_t> cls_of_;
};

// cudaMallocHost / cudaFreeHost replacements: pinned_take(&ptr, bytes),
// pinned_give(ptr)
template <typename T>
inline cudaError_t pinned_take(T **out, size_t bytes) {
  *out = static_cast<T *>(PinnedPool::get().take(bytes));
  return *out ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline void pinned_give(void *p) { PinnedPool::get().give(p); }

}  // namespace clgpu
