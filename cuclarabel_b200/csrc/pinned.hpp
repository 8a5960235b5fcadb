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
#include <cstdlib>
#include <iterator>
#include <map>
#include <mutex>
#include <new>
#include <utility>
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
        ++reused_;
        return p;
      }
    }
    void *p = nullptr;
    if (cudaMallocHost(&p, cls) != cudaSuccess) {
      cudaGetLastError();
      std::lock_guard<std::mutex> lk(mu_);
      ++failed_;
      return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu_);
    cls_of_[p] = cls;
    ++pinned_;
    pinned_bytes_ += (long long)cls;
    return p;
  }
  // takes served from the pool, page-locked allocations made, bytes
  // page-locked in all, failed allocations
  void stats(long long out[4]) {
    std::lock_guard<std::mutex> lk(mu_);
    out[0] = reused_;
    out[1] = pinned_;
    out[2] = pinned_bytes_;
    out[3] = failed_;
  }
  // returns p to the pool (false when p is not a pool buffer); a buffer
  // held for an owner's copies waits until the owner settles
  bool give(void *p) {
    if (!p) return false;
    std::lock_guard<std::mutex> lk(mu_);
    auto it = cls_of_.find(p);
    if (it == cls_of_.end()) return false;
    auto h = held_.find(p);
    if (h != held_.end()) {
      deferred_[h->second].push_back({p, it->second});
      held_.erase(h);
    } else {
      free_[it->second].push_back(p);
    }
    cls_of_.erase(it);
    return true;
  }
  bool owns(const void *p) {
    std::lock_guard<std::mutex> lk(mu_);
    return cls_of_.count(const_cast<void *>(p)) != 0;
  }
  // p (a pool buffer) is the source of asynchronous copies issued by
  // `owner`: if it is given back before the owner settles, it is kept out
  // of the pool until then
  void hold_for(void *p, const void *owner) {
    std::lock_guard<std::mutex> lk(mu_);
    if (cls_of_.count(p)) held_[p] = owner;
  }
  // the owner's copies have completed (its stream was synchronised)
  void settle(const void *owner) {
    std::lock_guard<std::mutex> lk(mu_);
    for (auto it = held_.begin(); it != held_.end();)
      it = it->second == owner ? held_.erase(it) : std::next(it);
    auto d = deferred_.find(owner);
    if (d == deferred_.end()) return;
    for (auto &e : d->second) free_[e.second].push_back(e.first);
    deferred_.erase(d);
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
  std::map<void *, const void *> held_;
  long long reused_ = 0, pinned_ = 0, pinned_bytes_ = 0, failed_ = 0;
  std::map<const void *, std::vector<std::pair<void *, size_t>>> deferred_;
};

// cudaMallocHost / cudaFreeHost replacements: pinned_take(&ptr, bytes),
// pinned_give(ptr)
template <typename T>
inline cudaError_t pinned_take(T **out, size_t bytes) {
  *out = static_cast<T *>(PinnedPool::get().take(bytes));
  return *out ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline void pinned_give(void *p) { PinnedPool::get().give(p); }

// Allocator of setup arrays: page-locked pool buffers (uploaded by
// asynchronous copies that overlap the rest of the setup), heap memory when
// no page-locked memory is left.  Elements are default-initialised (no zero
// fill): the arrays are written in full by parallel threads.
template <class T>
struct PinnedInitAlloc {
  using value_type = T;
  PinnedInitAlloc() = default;
  template <class U>
  PinnedInitAlloc(const PinnedInitAlloc<U> &) {}
  T *allocate(size_t n) {
    const size_t bytes = n * sizeof(T);
    void *p = PinnedPool::get().take(bytes);
    if (!p) p = std::malloc(bytes ? bytes : 1);
    if (!p) throw std::bad_alloc();
    return static_cast<T *>(p);
  }
  void deallocate(T *p, size_t) {
    if (!PinnedPool::get().give(p)) std::free(p);
  }
  template <class U>
  void construct(U *p) noexcept {
    ::new (static_cast<void *>(p)) U;
  }
  template <class U, class... Args>
  void construct(U *p, Args &&...args) {
    ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
  }
  template <class U>
  bool operator==(const PinnedInitAlloc<U> &) const {
    return true;
  }
  template <class U>
  bool operator!=(const PinnedInitAlloc<U> &) const {
    return false;
  }
};

}  // namespace clgpu
